"""Generate the golden fixtures in this folder from the reference's own code.

Runs only where the reference tree is present (the fixtures are committed, so
the tests never need it):
  1. unity_ell.json  -- the reference's unity/unity_ell.c, compiled from its
     sources by oracle/Makefile and run here: printed matrix, its, err, x.
     Also the same problem solved through the reference's ell_solve_jacobi via
     ctypes with every input initialised (b[9] = 0, x = 0), stored bit-exact.
  2. fem_tables.npz  -- the reference's fem_init tables (src/fem.c:61-408) and
     fem_init_struct 2D tables for two element sizes, read out of the
     reference's own globals.
  3. ell3d.npz       -- ELL matrices of small 3D meshes assembled with the
     reference's ell_init / ell_add_vals / ell_set_zero_row /
     ell_set_zero_col (src/ell.c) driven by the restated element loop of
     micro/src/assembly.c:93-135, and y = A x from the reference's ell_mvp
     for a seeded x (bit-exact).
  4. readme_2d.json  -- the 2D homogenized tensor printed in exs/README.md:
     154-157, with the run parameters.

    REF_DIR=<reference checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

# the reference checkout the fixtures are generated from (required)
REF_DIR = os.environ.get("REF_DIR", "")


def hexs(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def unity_ell():
    exe = O.REF_UNITY_ELL
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([exe], cwd=td, capture_output=True, text=True, check=True).stdout
        x_txt = open(os.path.join(td, "sol.dat")).read().split()
    lines = out.splitlines()
    i0 = lines.index("m=")
    mat = [[float(v) for v in ln.split()] for ln in lines[i0 + 1:i0 + 11]]
    its = int([ln for ln in lines if ln.startswith("its")][0].split("=")[1])
    err = float([ln for ln in lines if ln.startswith("err")][0].split("=")[1])
    # the same problem through the reference library with defined inputs
    R = O.ref()
    n = 10
    m = O.Ell()
    R.ell_init(C.byref(m), n, n, 4)
    me = np.array([1, -1, -1, 1], dtype=np.float64)
    b = np.zeros(n)
    for i in range(n - 1):
        b[i] = 1.0
        ix = np.array([i, i + 1], dtype=np.int32)
        R.ell_add_vals(C.byref(m), O.ptr(ix, O._ip), 2, O.ptr(ix, O._ip), 2, O.ptr(me))
    R.ell_set_zero_row(C.byref(m), 0, 1.0)
    R.ell_set_zero_row(C.byref(m), n - 1, 1.0)
    R.ell_set_zero_col(C.byref(m), 0, 1.0)
    R.ell_set_zero_col(C.byref(m), n - 1, 1.0)
    cols = np.ctypeslib.as_array(m.cols, shape=(n, 4)).copy()
    vals = np.ctypeslib.as_array(m.vals, shape=(n, 4)).copy()

    class Solver(C.Structure):
        _fields_ = [("max_its", C.c_int), ("its", C.c_int), ("min_err", C.c_double),
                    ("err", C.c_double)]

    R.ell_solve_jacobi.argtypes = [C.POINTER(Solver), C.POINTER(O.Ell), O._dp, O._dp]
    x = np.zeros(n)
    s = Solver()
    R.ell_solve_jacobi(C.byref(s), C.byref(m), O.ptr(b), O.ptr(x))
    return {
        "source": "unity/unity_ell.c run as compiled from the reference sources",
        "printed_matrix": mat, "printed_its": its, "printed_err": err,
        "printed_x": [float(v) for v in x_txt],
        "defined_inputs": {"b": hexs(b), "x0": hexs(np.zeros(n)), "its": s.its,
                           "err": float(s.err).hex(), "x": hexs(x),
                           "cols": cols.tolist(), "vals": hexs(vals)},
    }


def fem_tables():
    R = O.ref()
    R.fem_init.restype = C.c_int
    R.fem_init()
    out = {}
    dims = {"segm_2": (2, 1, 2), "tria_3": (3, 2, 3), "quad_4": (4, 2, 4), "tetra_4": (4, 3, 4),
            "prism_6": (6, 3, 6), "hexa_8": (8, 3, 8)}
    for name, (npe, dim, ngp) in dims.items():
        xp = C.POINTER(C.POINTER(C.c_double)).in_dll(R, f"xp_{name}")
        wp = C.POINTER(C.c_double).in_dll(R, f"wp_{name}")
        sh = C.POINTER(C.POINTER(C.c_double)).in_dll(R, f"sh_{name}")
        ds = C.POINTER(C.POINTER(C.POINTER(C.c_double))).in_dll(R, f"ds_{name}")
        out[f"xp_{name}"] = np.array([[xp[g][d] for d in range(dim)] for g in range(ngp)])
        out[f"wp_{name}"] = np.array([wp[g] for g in range(ngp)])
        out[f"sh_{name}"] = np.array([[sh[a][g] for g in range(ngp)] for a in range(npe)])
        out[f"ds_{name}"] = np.array([[[ds[a][d][g] for g in range(ngp)] for d in range(dim)]
                                      for a in range(npe)])
    R.fem_init_struct.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, O._dp, C.c_int]
    for tag, h in (("a", (0.25, 0.5)), ("b", (3.0 / 74, 3.0 / 74))):
        shp = C.POINTER(C.POINTER(C.c_double))()
        dshp = C.POINTER(C.POINTER(C.POINTER(C.c_double)))()
        wpp = C.POINTER(C.c_double)()
        hh = np.array(list(h) + [1.0])
        R.fem_init_struct(C.byref(shp), C.byref(dshp), C.byref(wpp), O.ptr(hh), 2)
        out[f"struct2d_{tag}_h"] = hh[:2]
        out[f"struct2d_{tag}_sh"] = np.array([[shp[a][g] for g in range(4)] for a in range(4)])
        out[f"struct2d_{tag}_dsh"] = np.array([[[dshp[a][d][g] for g in range(4)] for d in range(2)]
                                               for a in range(4)])
        out[f"struct2d_{tag}_wp"] = np.array([wpp[g] for g in range(4)])
    np.savez_compressed(os.path.join(HERE, "fem_tables.npz"), **out)


def ell3d():
    """Reference ELL assembly of small 3D meshes (n = 1, 2, 3 elements per edge)."""
    R = O.ref()
    out = {}
    E, nu = (1e9, 1e10), (0.3, 0.2)
    rng = np.random.default_rng(20261203)
    for n in (1, 2, 3):
        m = O.cube_mesh(n)
        et = O.fiber_types(m, [1.0, 1.0], 0.3 if n > 1 else 0.1)
        _, Ke, _, _ = O.operators(m, E, nu)
        A = O.Ell()
        R.ell_init(C.byref(A), m.ndof, m.ndof, 81)
        R.ell_set_zero_mat(C.byref(A))
        dofs = O.elem_dofs(m)
        for e in range(m.nelm):
            idx = np.ascontiguousarray(dofs[e])
            ke = np.ascontiguousarray(Ke[et[e]].reshape(-1))
            R.ell_add_vals(C.byref(A), O.ptr(idx, O._ip), 24, O.ptr(idx, O._ip), 24, O.ptr(ke))
        cols = np.ctypeslib.as_array(A.cols, shape=(m.ndof, 81)).copy()
        vals_raw = np.ctypeslib.as_array(A.vals, shape=(m.ndof, 81)).copy()
        # reference Dirichlet call sequence (micro/src/assembly.c:112-135, every boundary dof)
        for node in O.boundary_nodes(m):
            for d in range(3):
                R.ell_set_zero_row(C.byref(A), int(node) * 3 + d, 1.0)
                R.ell_set_zero_col(C.byref(A), int(node) * 3 + d, 1.0)
        vals_bc = np.ctypeslib.as_array(A.vals, shape=(m.ndof, 81)).copy()
        x = rng.standard_normal(m.ndof)
        y = np.zeros(m.ndof)
        R.ell_mvp(C.byref(A), O.ptr(x), O.ptr(y))
        out[f"n{n}_etype"] = et
        out[f"n{n}_cols"] = cols
        out[f"n{n}_vals_raw"] = vals_raw
        out[f"n{n}_vals_bc"] = vals_bc
        out[f"n{n}_x"] = x
        out[f"n{n}_y"] = y
    np.savez_compressed(os.path.join(HERE, "ell3d.npz"), **out)


def readme_2d():
    return {
        "source": "exs/README.md:136-157 (micro_alone example, printed tensor)",
        "struct_n_nodes": [75, 75], "size": [3.0, 3.0],
        "materials": {"MATRIX": {"rho": 1e7, "E": 1e6, "nu": 0.3},
                      "FIBER": {"rho": 1e7, "E": 1e7, "nu": 0.3}},
        "command_line_radius": 0.75,
        "reproducing_radius": 0.9,
        "C": [[2.050980e+06, 7.787895e+05, 0.0], [7.786073e+05, 2.050987e+06, 0.0],
              [0.0, 0.0, 6.080510e+05]],
        "note": ("printed with %e (7 significant digits) after a PETSc CG solve of unknown "
                 "tolerance; the current code reproduces it with radius 0.9, not the 0.75 "
                 "of the printed command line"),
    }


def main():
    if not REF_DIR or not os.path.isdir(REF_DIR):
        sys.exit("set REF_DIR to the reference checkout (the fixtures are committed)")
    os.environ["REF_DIR"] = REF_DIR
    O.build()
    json.dump(unity_ell(), open(os.path.join(HERE, "unity_ell.json"), "w"), indent=1)
    fem_tables()
    ell3d()
    json.dump(readme_2d(), open(os.path.join(HERE, "readme_2d.json"), "w"), indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()

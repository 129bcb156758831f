"""ctypes binding of the CPU oracle (oracle.c) and of the reference's own
ell.c / fem.c compiled from its sources (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker or the timed CPU baseline.  The
product library (madmax_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref.so")
REF_UNITY_ELL = os.path.join(HERE, "_ref", "unity_ell")

ID_MATRIX, ID_FIBER = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_ubyte)


class Mesh(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "dim", "nx", "ny", "nz", "nex", "ney", "nez", "nelm", "nn", "npe", "nvoi", "ngp", "ndof")
    ] + [(n, C.c_double) for n in ("lx", "ly", "lz", "hx", "hy", "hz", "vol", "vol_elm")]


class Ell(C.Structure):
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("nnz", C.c_int),
                ("cols", _ip), ("vals", _dp)]


class Params(C.Structure):
    _fields_ = [("E", C.c_double * 2), ("nu", C.c_double * 2), ("rtol", C.c_double),
                ("lin_rtol", C.c_double), ("max_newton", C.c_int), ("max_lin_its", C.c_int),
                ("solver", C.c_int)]


def build(force: bool = False) -> None:
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    args = ["make", "-s", "-C", HERE] + (["-B"] if force else [])
    subprocess.run(args, check=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_mesh_init.argtypes = [C.POINTER(Mesh), C.c_int, _ip, _dp]
        L.orc_elem_dofs.argtypes = [C.POINTER(Mesh), C.c_int, _ip]
        L.orc_elem_nodes.argtypes = [C.POINTER(Mesh), C.c_int, _ip]
        L.orc_is_boundary_node.argtypes = [C.POINTER(Mesh), C.c_int]
        L.orc_boundary_nodes.argtypes = [C.POINTER(Mesh), _ip]
        L.orc_fiber_cilin_types.argtypes = [C.POINTER(Mesh), _dp, C.c_int, C.c_int, C.c_double,
                                            _dp, _up]
        L.orc_hexa8_tables.argtypes = [_dp, _dp, _dp]
        L.orc_struct_dsh.argtypes = [C.POINTER(Mesh), _dp, _dp]
        L.orc_bmat.argtypes = [C.POINTER(Mesh), _dp, _dp]
        L.orc_iso_D.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
        L.orc_elem_stiffness.argtypes = [C.POINTER(Mesh), _dp, _dp, _dp, _dp]
        L.orc_ell_init.argtypes = [C.POINTER(Ell), C.c_int, C.c_int, C.c_int]
        L.orc_ell_free.argtypes = [C.POINTER(Ell)]
        L.orc_ell_mvp.argtypes = [C.POINTER(Ell), _dp, _dp]
        L.orc_assemble_jac.argtypes = [C.POINTER(Mesh), _up, _dp, C.POINTER(Ell), C.c_int]
        L.orc_assemble_res.argtypes = [C.POINTER(Mesh), _up, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_affine_bc.argtypes = [C.POINTER(Mesh), _dp, _dp]
        L.orc_averages.argtypes = [C.POINTER(Mesh), _up, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_jacobi.argtypes = [C.POINTER(Ell), _dp, _dp, C.c_int, C.c_double, _ip, _dp]
        L.orc_pcg.argtypes = [C.POINTER(Ell), _dp, _dp, C.c_double, C.c_int, _ip, _dp]
        L.orc_homogenize.argtypes = [C.POINTER(Mesh), _up, C.POINTER(Params), C.c_int, _dp, _dp,
                                     _dp, _dp, _dp]
        L.orc_unit_tangent.argtypes = [C.POINTER(Mesh), _up, C.POINTER(Params), _dp, _dp]
        L.orc_fd_tangent.argtypes = [C.POINTER(Mesh), _up, C.POINTER(Params), _dp, _dp, _dp]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref():
    """The reference's own ell.c/fem.c (compiled unchanged)."""
    global _ref
    if _ref is None:
        R = C.CDLL(REF_LIB_PATH)
        R.ell_init.argtypes = [C.POINTER(Ell), C.c_int, C.c_int, C.c_int]
        R.ell_add_vals.argtypes = [C.POINTER(Ell), _ip, C.c_int, _ip, C.c_int, _dp]
        R.ell_set_zero_row.argtypes = [C.POINTER(Ell), C.c_int, C.c_double]
        R.ell_set_zero_col.argtypes = [C.POINTER(Ell), C.c_int, C.c_double]
        R.ell_set_zero_mat.argtypes = [C.POINTER(Ell)]
        R.ell_mvp.argtypes = [C.POINTER(Ell), _dp, _dp]
        R.ell_get_val.argtypes = [C.POINTER(Ell), C.c_int, C.c_int, _dp]
        _ref = R
    return _ref


def ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------- helpers ---

def mesh(dim: int, n_nodes, length) -> Mesh:
    m = Mesh()
    nn = np.ascontiguousarray(n_nodes, dtype=np.int32)
    ln = np.ascontiguousarray(length, dtype=np.float64)
    rc = lib().orc_mesh_init(C.byref(m), dim, ptr(nn, _ip), ptr(ln))
    if rc:
        raise ValueError(f"orc_mesh_init failed ({rc})")
    return m


def cube_mesh(n: int, length: float = 1.0) -> Mesh:
    """3D unit cube with n elements per edge (n+1 nodes)."""
    return mesh(3, [n + 1] * 3, [length] * 3)


def fiber_types(m: Mesh, size, radius: float, nfib=(1, 1), desv=(0.0, 0.0)) -> np.ndarray:
    et = np.zeros(m.nelm, dtype=np.uint8)
    sz = np.ascontiguousarray(size, dtype=np.float64)
    dv = np.ascontiguousarray(desv, dtype=np.float64)
    lib().orc_fiber_cilin_types(C.byref(m), ptr(sz), nfib[0], nfib[1], radius, ptr(dv),
                                ptr(et, _up))
    return et


def elem_dofs(m: Mesh) -> np.ndarray:
    nc = m.npe * m.dim
    out = np.zeros((m.nelm, nc), dtype=np.int32)
    tmp = np.zeros(nc, dtype=np.int32)
    for e in range(m.nelm):
        lib().orc_elem_dofs(C.byref(m), e, ptr(tmp, _ip))
        out[e] = tmp
    return out


def boundary_nodes(m: Mesh) -> np.ndarray:
    c = lib().orc_boundary_nodes(C.byref(m), None)
    out = np.zeros(c, dtype=np.int32)
    lib().orc_boundary_nodes(C.byref(m), ptr(out, _ip))
    return out


def operators(m: Mesh, E, nu):
    """(D_by_type [2,nvoi,nvoi], Ke_by_type [2,nc,nc], bmat, wp)."""
    nvoi, nc, ngp = m.nvoi, m.npe * m.dim, m.ngp
    dsh = np.zeros(m.npe * m.dim * ngp)
    wp = np.zeros(ngp)
    lib().orc_struct_dsh(C.byref(m), ptr(dsh), ptr(wp))
    bmat = np.zeros(nvoi * nc * ngp)
    lib().orc_bmat(C.byref(m), ptr(dsh), ptr(bmat))
    D = np.zeros((2, nvoi * nvoi))
    Ke = np.zeros((2, nc * nc))
    for t in range(2):
        Dt = np.zeros(nvoi * nvoi)
        lib().orc_iso_D(m.dim, E[t], nu[t], ptr(Dt))
        D[t] = Dt
        Kt = np.zeros(nc * nc)
        lib().orc_elem_stiffness(C.byref(m), ptr(bmat), ptr(wp), ptr(Dt), ptr(Kt))
        Ke[t] = Kt
    return D.reshape(2, nvoi, nvoi), Ke.reshape(2, nc, nc), bmat, wp


class EllMatrix:
    """Owning wrapper around an orc_ell."""

    def __init__(self, nrow, ncol, width):
        self.s = Ell()
        if lib().orc_ell_init(C.byref(self.s), nrow, ncol, width):
            raise MemoryError("orc_ell_init")
        self.nrow, self.width = nrow, width

    @property
    def cols(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.s.cols, shape=(self.nrow, self.width))

    @property
    def vals(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.s.vals, shape=(self.nrow, self.width))

    def mvp(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.nrow)
        lib().orc_ell_mvp(C.byref(self.s), ptr(x), ptr(y))
        return y

    def __del__(self):
        try:
            lib().orc_ell_free(C.byref(self.s))
        except Exception:
            pass


def assemble(m: Mesh, etype: np.ndarray, E, nu, symmetric_bc: bool = True) -> EllMatrix:
    _, Ke, _, _ = operators(m, E, nu)
    width = 18 if m.dim == 2 else 81
    A = EllMatrix(m.ndof, m.ndof, width)
    Kf = np.ascontiguousarray(Ke.reshape(-1))
    lib().orc_assemble_jac(C.byref(m), ptr(etype, _up), ptr(Kf), C.byref(A.s), int(symmetric_bc))
    return A


def affine_bc(m: Mesh, strain) -> np.ndarray:
    u = np.zeros(m.ndof)
    s = np.ascontiguousarray(strain, dtype=np.float64)
    lib().orc_affine_bc(C.byref(m), ptr(s), ptr(u))
    return u


def residual(m: Mesh, etype, E, nu, u):
    D, _, bmat, wp = operators(m, E, nu)
    Df = np.ascontiguousarray(D.reshape(-1))
    r = np.zeros(m.ndof)
    nrm = C.c_double()
    lib().orc_assemble_res(C.byref(m), ptr(etype, _up), ptr(Df), ptr(bmat), ptr(wp),
                           ptr(np.ascontiguousarray(u, dtype=np.float64)), ptr(r), C.byref(nrm))
    return r, nrm.value


def averages(m: Mesh, etype, E, nu, u):
    D, _, bmat, wp = operators(m, E, nu)
    Df = np.ascontiguousarray(D.reshape(-1))
    sa = np.zeros(m.nvoi)
    st = np.zeros(m.nvoi)
    lib().orc_averages(C.byref(m), ptr(etype, _up), ptr(Df), ptr(bmat), ptr(wp),
                       ptr(np.ascontiguousarray(u, dtype=np.float64)), ptr(sa), ptr(st))
    return sa, st


def params(E, nu, rtol=1e-8, lin_rtol=1e-9, max_newton=4, max_lin_its=100000, solver=0) -> Params:
    p = Params()
    p.E[0], p.E[1] = E
    p.nu[0], p.nu[1] = nu
    p.rtol, p.lin_rtol = rtol, lin_rtol
    p.max_newton, p.max_lin_its, p.solver = max_newton, max_lin_its, solver
    return p


def homogenize(m: Mesh, etype, E, nu, strains, want_u=False, **kw):
    """Returns (strain_ave [k,nvoi], stress_ave [k,nvoi], u [k,ndof] | None, stats [k,4])."""
    strains = np.ascontiguousarray(np.atleast_2d(strains), dtype=np.float64)
    k = strains.shape[0]
    sa = np.zeros((k, m.nvoi))
    st = np.zeros((k, m.nvoi))
    stats = np.zeros((k, 4))
    u = np.zeros((k, m.ndof)) if want_u else None
    p = params(E, nu, **kw)
    rc = lib().orc_homogenize(C.byref(m), ptr(etype, _up), C.byref(p), k, ptr(strains), ptr(sa),
                              ptr(st), ptr(u) if want_u else None, ptr(stats))
    if rc:
        raise RuntimeError(f"orc_homogenize failed ({rc})")
    return sa, st, u, stats


def unit_tangent(m: Mesh, etype, E, nu, **kw):
    C6 = np.zeros(m.nvoi * m.nvoi)
    stats = np.zeros(m.nvoi * 4)
    p = params(E, nu, **kw)
    rc = lib().orc_unit_tangent(C.byref(m), ptr(etype, _up), C.byref(p), ptr(C6), ptr(stats))
    if rc:
        raise RuntimeError(f"orc_unit_tangent failed ({rc})")
    return C6.reshape(m.nvoi, m.nvoi), stats.reshape(m.nvoi, 4)


def fd_tangent(m: Mesh, etype, E, nu, strain_mac, **kw):
    C6 = np.zeros(m.nvoi * m.nvoi)
    s0 = np.zeros(m.nvoi)
    p = params(E, nu, **kw)
    sm = np.ascontiguousarray(strain_mac, dtype=np.float64)
    rc = lib().orc_fd_tangent(C.byref(m), ptr(etype, _up), C.byref(p), ptr(sm), ptr(C6), ptr(s0))
    if rc:
        raise RuntimeError(f"orc_fd_tangent failed ({rc})")
    return C6.reshape(m.nvoi, m.nvoi), s0

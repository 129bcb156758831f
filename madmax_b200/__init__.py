"""madmax_b200 -- Python view of libsputnik_b200.so, the B200 (sm_100a)
implementation of sputnik's micro-RVE homogenization hot path.

The product is the C ABI in include/*.h; this module binds it with ctypes for
the tests, the benchmark and Python callers.  It has no compute of its own and
no fallback: if the shared library is missing it raises at import, and without
a CUDA device the compute calls raise SputnikError(SP_ERR_CUDA).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsputnik_b200.so")

SP_OK, SP_ERR_ARG, SP_ERR_NOMEM, SP_ERR_RANGE = 0, 1, 2, 3
SP_ERR_CUDA, SP_ERR_NOCONV, SP_ERR_BUDGET, SP_ERR_TIMEOUT, SP_ERR_STATE, SP_PENDING = 5, 6, 7, 8, 9, 10
ELL_ERR_CUDA = 5
SP_ID_MATRIX, SP_ID_FIBER = 0, 1
SP_PREC_MIXED, SP_PREC_FP64 = 0, 1
SP_OP_ELL, SP_OP_STENCIL = 0, 1
SP_BC_AFFINE, SP_BC_PERIODIC = 0, 1
SP_TUNE_AUTO, SP_TUNE_OFF = 0, 1
SP_MAX_RHS = 8
SP_NOALLOC_MAX_ROWS = 262144
MAX_ITS, MIN_ERR = 100000, 1.0e-10

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_ubyte)
_vp = C.c_void_p


class SputnikError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


# ------------------------------------------------------------------ structs ---

class ell_matrix(C.Structure):
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("nnz", C.c_int), ("cols", _ip),
                ("vals", _dp)]


class ell_solver(C.Structure):
    _fields_ = [("max_its", C.c_int), ("its", C.c_int), ("min_err", C.c_double),
                ("err", C.c_double)]


class sp_rve_desc(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("len", C.c_double * 3), ("nx_fib", C.c_int),
                ("ny_fib", C.c_int), ("radius", C.c_double), ("desv", C.c_double * 2),
                ("E", C.c_double * 2), ("nu", C.c_double * 2)]


class sp_solve_info(C.Structure):
    _fields_ = [("status", C.c_int), ("outer_its", C.c_int), ("inner_its", C.c_int),
                ("pad", C.c_int), ("relres", C.c_double)]


class sp_batch_opts(C.Structure):
    _fields_ = [("nrhs", C.c_int), ("precision", C.c_int), ("rtol", C.c_double),
                ("inner_rtol", C.c_double), ("max_outer", C.c_int), ("max_inner", C.c_int),
                ("threads", C.c_int), ("lanes_per_row", C.c_int), ("ctas_per_sm", C.c_int),
                ("cluster", C.c_int), ("op", C.c_int), ("bc", C.c_int), ("tune", C.c_int)]


class sp_server_opts(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_inflight", C.c_int),
                ("queue_capacity", C.c_int), ("rtol", C.c_double), ("inner_rtol", C.c_double),
                ("idle_spin_limit", C.c_int), ("op", C.c_int), ("ctas_per_sm", C.c_int),
                ("refine_rtol", C.c_double), ("warm_start", C.c_int)]


SP_ACTION_NULL, SP_ACTION_MICRO_CALC_STRESS, SP_ACTION_MICRO_CALC_C_TANGENT = 0, 1, 2
SP_ACTION_MICRO_CALC_RHO, SP_ACTION_MICRO_END = 3, 4
SP_MICRO_LINEAR, SP_MICRO_SOLVE = 0, 1
SP_WARM_PREDICT, SP_WARM_LAST = 0, 1


class sp_message(C.Structure):
    """message_t of the reference (inc/comm.h:18-27)."""
    _fields_ = [("action", C.c_int), ("num_voigt", C.c_int), ("strain_mac", C.c_double * 6),
                ("stress_ave", C.c_double * 6), ("c_tangent_ave", C.c_double * 36),
                ("rho", C.c_double)]


MESSAGE_RECV = C.CFUNCTYPE(C.c_int, C.POINTER(sp_message), C.c_void_p)
MESSAGE_SEND = C.CFUNCTYPE(C.c_int, C.POINTER(sp_message), C.c_void_p)

SP_FE2_LINEAR, SP_FE2_PER_GP, SP_FE2_MAX_ITS = 0, 1, 16


class sp_fe2_desc(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("len", C.c_double * 3), ("traction", C.c_double * 3),
                ("nrve", C.c_int), ("rves", C.POINTER(sp_rve_desc)), ("gp_rve", C.POINTER(C.c_int)),
                ("newton_its", C.c_int), ("newton_tol", C.c_double), ("lin_rtol", C.c_double),
                ("strain_clip", C.c_double), ("micro", C.c_int), ("seed", C.c_int)]


class sp_fe2_info(C.Structure):
    _fields_ = [("newton_its", C.c_int), ("pcg_its", C.c_int * 16), ("bnorm", C.c_double * 16),
                ("tip", C.c_double * 3), ("micro_requests", C.c_longlong),
                ("micro_s", C.c_double), ("macro_s", C.c_double), ("residual_ms", C.c_double),
                ("assemble_ms", C.c_double), ("solve_ms", C.c_double)]


# ------------------------------------------------------------------- loader ---

# name -> (restype, argtypes); every symbol the public headers declare
_PROTOS = {
    # ell.h
    "ell_init": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_int, C.c_int]),
    "ell_set_val": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_int, C.c_double]),
    "ell_add_val": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_int, C.c_double]),
    "ell_add_vals": (C.c_int, [C.POINTER(ell_matrix), _ip, C.c_int, _ip, C.c_int, _dp]),
    "ell_mvp": (C.c_int, [C.POINTER(ell_matrix), _dp, _dp]),
    "ell_get_val": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_int, _dp]),
    "ell_solve_jacobi": (C.c_int, [C.POINTER(ell_solver), C.POINTER(ell_matrix), _dp, _dp]),
    "ell_set_zero_row": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_double]),
    "ell_set_zero_col": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_double]),
    "ell_set_zero_mat": (C.c_int, [C.POINTER(ell_matrix)]),
    "ell_print_full": (C.c_int, [C.POINTER(ell_matrix)]),
    # fem.h
    "fem_init": (C.c_int, []),
    "fem_init_struct": (C.c_int, [_vp, _vp, _vp, _dp, C.c_int]),
    "fem_invjac": (C.c_int, [C.c_int, _vp, _vp, _dp]),
    "fem_calc_jac": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _vp, _vp]),
    "fem_trans_dsh": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "fem_get_dsh_master": (C.c_int, [C.c_int, C.c_int, _vp]),
    "fem_get_sh": (C.c_int, [C.c_int, C.c_int, _vp]),
    "fem_get_wp": (C.c_int, [C.c_int, C.c_int, _vp]),
    # sputnik_b200.h
    "sp_last_error": (C.c_char_p, []),
    "sp_version": (C.c_int, []),
    "sp_init": (C.c_int, [C.c_int]),
    "sp_device_count": (C.c_int, []),
    "ell_set_zero_col_full": (C.c_int, [C.POINTER(ell_matrix), C.c_int, C.c_double]),
    "ell_free": (C.c_int, [C.POINTER(ell_matrix)]),
    "sp_ell_upload": (C.c_int, [C.POINTER(ell_matrix), C.POINTER(_vp)]),
    "sp_ell_dev_free": (C.c_int, [_vp]),
    "sp_ell_dev_mvp": (C.c_int, [_vp, _vp, _vp, _vp]),
    "sp_ell_dev_mvp_host": (C.c_int, [_vp, _dp, _dp]),
    "sp_ell_dev_set_lanes": (C.c_int, [_vp, C.c_int]),
    "sp_ell_dev_info": (C.c_int, [_vp, _ip, _ip, C.POINTER(C.c_longlong)]),
    "sp_ell_dev_pcg": (C.c_int, [_vp, _dp, _dp, C.c_double, C.c_int, _ip, _dp]),
    "sp_ell_pcg_noalloc": (C.c_int, [C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_double, C.c_int,
                                     _ip, _dp, _vp]),
    "sp_classify": (C.c_int, [C.POINTER(sp_rve_desc), _up]),
    "sp_rve_fields": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp]),
    "sp_micro_create": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.POINTER(_vp)]),
    "sp_micro_destroy": (C.c_int, [_vp]),
    "sp_micro_handle": (C.c_int, [_vp, C.POINTER(sp_message)]),
    "sp_micro_serve": (C.c_int, [_vp, MESSAGE_RECV, MESSAGE_SEND, C.c_void_p,
                                 C.POINTER(C.c_longlong)]),
    "sp_micro_requests": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "sp_rve_write_vtu": (C.c_int, [_vp, C.c_int, C.c_char_p]),
    "sp_vtu_write": (C.c_int, [C.c_char_p, _ip, _dp, _dp, _dp, _up, _dp, _dp]),
    "sp_fe2_desc_default": (None, [C.POINTER(sp_fe2_desc)]),
    "sp_fe2_create": (C.c_int, [C.POINTER(sp_fe2_desc), C.POINTER(_vp)]),
    "sp_fe2_run": (C.c_int, [_vp, C.POINTER(sp_fe2_info)]),
    "sp_fe2_displacement": (C.c_int, [_vp, _dp]),
    "sp_fe2_gp_rve": (C.c_int, [_vp, _ip]),
    "sp_fe2_micro_tangents": (C.c_int, [_vp, _dp]),
    "sp_fe2_destroy": (C.c_int, [_vp]),
    "sp_ell_pattern": (C.c_int, [_ip, _ip]),
    "sp_rve_create": (C.c_int, [C.POINTER(sp_rve_desc), C.POINTER(_vp)]),
    "sp_rve_destroy": (C.c_int, [_vp]),
    "sp_rve_sizes": (C.c_int, [_vp, _ip, _ip, _ip]),
    "sp_rve_get_ell": (C.c_int, [_vp, _ip, _dp]),
    "sp_rve_get_ke": (C.c_int, [_vp, _dp, _dp]),
    "sp_rve_homogenize": (C.c_int, [_vp, C.c_int, _dp, C.c_double, _dp, _dp, _dp,
                                    C.POINTER(sp_solve_info)]),
    "sp_rve_tangent": (C.c_int, [_vp, C.c_double, _dp, C.POINTER(sp_solve_info)]),
    "sp_batch_opts_default": (None, [C.POINTER(sp_batch_opts)]),
    "sp_batch_create": (C.c_int, [C.c_int, C.POINTER(sp_rve_desc), C.POINTER(sp_batch_opts),
                                  C.POINTER(_vp)]),
    "sp_batch_destroy": (C.c_int, [_vp]),
    "sp_batch_set_etype": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_ubyte), _vp]),
    "sp_batch_device_bytes": (C.c_int, [_vp, C.POINTER(C.c_size_t)]),
    "sp_batch_shape": (C.c_int, [_vp, _ip, _ip, _ip]),
    "sp_batch_tune_report": (C.c_int, [_vp, C.c_int, _ip, _ip, _dp, _ip, _ip, _ip]),
    "sp_ell_dev_lanes": (C.c_int, [_vp, _ip, C.POINTER(C.c_float), _ip]),
    "sp_server_status": (C.c_int, [_vp, _ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sp_batch_upload": (C.c_int, [_vp, _dp, _dp, _vp]),
    "sp_batch_launch": (C.c_int, [_vp, _vp]),
    "sp_batch_download": (C.c_int, [_vp, _dp, _dp, C.POINTER(sp_solve_info), _vp]),
    "sp_batch_homogenize": (C.c_int, [_vp, _dp, _dp, _dp, _dp, C.POINTER(sp_solve_info), _vp]),
    "sp_batch_last_launches": (C.c_int, [_vp, _ip]),
    "sp_server_opts_default": (None, [C.POINTER(sp_server_opts)]),
    "sp_server_create": (C.c_int, [C.c_int, C.POINTER(sp_rve_desc), C.POINTER(sp_server_opts),
                                   C.POINTER(_vp)]),
    "sp_server_destroy": (C.c_int, [_vp]),
    "sp_server_plan_bytes": (C.c_int, [C.c_int, C.POINTER(sp_rve_desc),
                                       C.POINTER(sp_server_opts), C.POINTER(C.c_size_t)]),
    "sp_server_start": (C.c_int, [_vp]),
    "sp_server_submit": (C.c_int, [_vp, C.c_int, _dp, C.POINTER(C.c_longlong)]),
    "sp_server_poll": (C.c_int, [_vp, C.c_longlong, _dp, _dp, C.POINTER(sp_solve_info)]),
    "sp_server_stop": (C.c_int, [_vp]),
    "sp_server_replay": (C.c_int, [_vp, C.c_int, _ip, _dp, _dp, _dp, _dp, _dp,
                                   C.POINTER(sp_solve_info), C.c_double]),
}

# data symbols the headers declare (fem.h tables, solvers.h selector)
DATA_SYMBOLS = [f"{k}_{e}" for e in ("segm_2", "tria_3", "quad_4", "tetra_4", "prism_6", "hexa_8")
                for k in ("xp", "wp", "sh", "ds")] + ["solver"]

_lib = None
MISSING: list = []  # prototypes the loaded library does not export


def load() -> C.CDLL:
    """Load libsputnik_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run `python -m madmax_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            try:
                f = getattr(L, name)
            except AttributeError:
                MISSING.append(name)
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def lib() -> C.CDLL:
    return load()


def last_error() -> str:
    return (lib().sp_last_error() or b"").decode()


def check(rc: int, what: str = "") -> None:
    if rc != 0 and rc != SP_PENDING:
        raise SputnikError(rc, f"{what}: {last_error()}")


def device_count() -> int:
    return lib().sp_device_count()


def ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


# --------------------------------------------------------------- ELL (drop-in)

class EllMatrix:
    """Owns an ell_matrix built by the library's ell_init (host arrays)."""

    def __init__(self, nrow: int, ncol: int, nnz: int):
        self.m = ell_matrix()
        check(lib().ell_init(C.byref(self.m), nrow, ncol, nnz), "ell_init")

    @property
    def cols(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.m.cols, shape=(self.m.nrow, self.m.nnz))

    @property
    def vals(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.m.vals, shape=(self.m.nrow, self.m.nnz))

    def add_vals(self, ix, iy, vals) -> int:
        ix = np.ascontiguousarray(ix, dtype=np.int32)
        iy = np.ascontiguousarray(iy, dtype=np.int32)
        v = np.ascontiguousarray(vals, dtype=np.float64)
        return lib().ell_add_vals(C.byref(self.m), ptr(ix, _ip), len(ix), ptr(iy, _ip), len(iy),
                                  ptr(v))

    def mvp(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.m.nrow)
        check(lib().ell_mvp(C.byref(self.m), ptr(x), ptr(y)), "ell_mvp")
        return y

    def solve_jacobi(self, b, x0):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64)
        s = ell_solver()
        check(lib().ell_solve_jacobi(C.byref(s), C.byref(self.m), ptr(b), ptr(x)),
              "ell_solve_jacobi")
        return x, s.its, s.err

    def __del__(self):
        try:
            lib().ell_free(C.byref(self.m))
        except Exception:
            pass


# ---------------------------------------------------------------------- RVE

def rve_desc(n, radius=0.25, E=(1e9, 1e10), nu=(0.3, 0.2), length=1.0, nfib=(1, 1),
             desv=(0.0, 0.0)) -> sp_rve_desc:
    d = sp_rve_desc()
    nn = (n, n, n) if np.isscalar(n) else tuple(n)
    ll = (length,) * 3 if np.isscalar(length) else tuple(length)
    for k in range(3):
        d.n[k] = int(nn[k])
        d.len[k] = float(ll[k])
    d.nx_fib, d.ny_fib = nfib
    d.radius = radius
    d.desv[0], d.desv[1] = desv
    d.E[0], d.E[1] = E
    d.nu[0], d.nu[1] = nu
    return d


def classify(desc: sp_rve_desc) -> np.ndarray:
    nelm = desc.n[0] * desc.n[1] * desc.n[2]
    et = np.zeros(nelm, dtype=np.uint8)
    check(lib().sp_classify(C.byref(desc), ptr(et, _up)), "sp_classify")
    return et


def ell_pattern(n) -> np.ndarray:
    nn = np.array([n] * 3 if np.isscalar(n) else n, dtype=np.int32)
    ndof = 3 * int(np.prod(nn + 1))
    cols = np.zeros((ndof, 81), dtype=np.int32)
    check(lib().sp_ell_pattern(ptr(nn, _ip), ptr(cols, _ip)), "sp_ell_pattern")
    return cols


class Rve:
    """One RVE on the GPU (plain FP64 path)."""

    def __init__(self, desc: sp_rve_desc):
        self.desc = desc
        self.h = _vp()
        check(lib().sp_rve_create(C.byref(desc), C.byref(self.h)), "sp_rve_create")
        nd, ne, nf = C.c_int(), C.c_int(), C.c_int()
        check(lib().sp_rve_sizes(self.h, C.byref(nd), C.byref(ne), C.byref(nf)), "sp_rve_sizes")
        self.ndof, self.nelm, self.nfiber = nd.value, ne.value, nf.value

    def ell(self):
        cols = np.zeros((self.ndof, 81), dtype=np.int32)
        vals = np.zeros((self.ndof, 81))
        check(lib().sp_rve_get_ell(self.h, ptr(cols, _ip), ptr(vals)), "sp_rve_get_ell")
        return cols, vals

    def ke(self):
        a = np.zeros(576)
        b = np.zeros(576)
        check(lib().sp_rve_get_ke(self.h, ptr(a), ptr(b)), "sp_rve_get_ke")
        return a.reshape(24, 24), b.reshape(24, 24)

    def homogenize(self, strains, rtol=1e-8, want_u=False):
        s = np.ascontiguousarray(np.atleast_2d(strains), dtype=np.float64)
        k = s.shape[0]
        sa = np.zeros((k, 6))
        st = np.zeros((k, 6))
        u = np.zeros((k, self.ndof)) if want_u else None
        info = sp_solve_info()
        check(lib().sp_rve_homogenize(self.h, k, ptr(s), rtol, ptr(sa), ptr(st), ptr(u),
                                      C.byref(info)), "sp_rve_homogenize")
        return sa, st, u, info

    def tangent(self, rtol=1e-8):
        Cm = np.zeros(36)
        info = sp_solve_info()
        check(lib().sp_rve_tangent(self.h, rtol, ptr(Cm), C.byref(info)), "sp_rve_tangent")
        return Cm.reshape(6, 6), info

    def fields(self, q=0):
        """(strain_e [nelm,6], stress_e [nelm,6], u [ndof], residual [ndof]) of
        load case q of the last solve."""
        se, st = np.zeros((self.nelm, 6)), np.zeros((self.nelm, 6))
        u, r = np.zeros(self.ndof), np.zeros(self.ndof)
        check(lib().sp_rve_fields(self.h, q, ptr(se), ptr(st), ptr(u), ptr(r)), "sp_rve_fields")
        return se, st, u, r

    def write_vtu(self, base: str, q=0):
        check(lib().sp_rve_write_vtu(self.h, q, base.encode()), "sp_rve_write_vtu")

    def close(self):
        if self.h:
            lib().sp_rve_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -------------------------------------------------------------------- batch

def batch_opts(**kw) -> sp_batch_opts:
    o = sp_batch_opts()
    lib().sp_batch_opts_default(C.byref(o))
    names = {f[0] for f in sp_batch_opts._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError(f"unknown batch option {k!r}")
        setattr(o, k, v)
    return o


class Batch:
    """Many RVEs solved by one persistent launch (mixed precision by default)."""

    def __init__(self, descs, **opts):
        self.n = len(descs)
        self.descs = (sp_rve_desc * self.n)(*descs)
        self.opts = batch_opts(**opts)
        self.h = _vp()
        check(lib().sp_batch_create(self.n, self.descs, C.byref(self.opts), C.byref(self.h)),
              "sp_batch_create")
        self.nrhs = self.opts.nrhs

    def shape(self):
        """(threads per CTA, CTAs per SM, persistent grid)."""
        t, c, g = C.c_int(), C.c_int(), C.c_int()
        check(lib().sp_batch_shape(self.h, C.byref(t), C.byref(c), C.byref(g)), "sp_batch_shape")
        return t.value, c.value, g.value

    def tune_report(self) -> dict:
        """The autotuner's trial: candidate shapes with their measured rates
        (estimated work units per ms), the chosen one, and whether it came
        from the process-wide cache; empty when the shape was given."""
        th = (C.c_int * 8)()
        ct = (C.c_int * 8)()
        rt = (C.c_double * 8)()
        n, ch, fc = C.c_int(), C.c_int(), C.c_int()
        check(lib().sp_batch_tune_report(self.h, 8, th, ct, rt, C.byref(n), C.byref(ch),
                                         C.byref(fc)), "sp_batch_tune_report")
        if n.value == 0:
            return {}
        return {"candidates": [{"threads": th[k], "ctas_per_sm": ct[k], "rate": rt[k]}
                               for k in range(n.value)],
                "chosen": {"threads": th[ch.value], "ctas_per_sm": ct[ch.value]},
                "from_cache": bool(fc.value)}

    def device_bytes(self) -> int:
        b = C.c_size_t()
        check(lib().sp_batch_device_bytes(self.h, C.byref(b)), "sp_batch_device_bytes")
        return b.value

    def upload(self, strains=None, materials=None, stream=None):
        check(lib().sp_batch_upload(self.h, ptr(strains), ptr(materials), stream),
              "sp_batch_upload")

    def set_etype(self, rve: int, etype, stream=None):
        """Element materials of RVE `rve` (0 matrix, 1 fibre, x-fastest) in
        place of its fibre classification, from the next launch on."""
        et = np.ascontiguousarray(etype, dtype=np.uint8)
        check(lib().sp_batch_set_etype(self.h, int(rve), et.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                       stream), "sp_batch_set_etype")

    def launch(self, stream=None):
        check(lib().sp_batch_launch(self.h, stream), "sp_batch_launch")

    def download(self, stress=None, strain=None, info=None, stream=None):
        check(lib().sp_batch_download(self.h, ptr(stress), ptr(strain), info, stream),
              "sp_batch_download")

    def homogenize(self, strains=None, materials=None, stream=None):
        stress = np.zeros((self.n, self.nrhs, 6))
        strain = np.zeros((self.n, self.nrhs, 6))
        info = (sp_solve_info * self.n)()
        check(lib().sp_batch_homogenize(self.h, ptr(strains), ptr(materials), ptr(stress),
                                        ptr(strain), info, stream), "sp_batch_homogenize")
        return stress, strain, info

    def last_launches(self) -> int:
        n = C.c_int()
        check(lib().sp_batch_last_launches(self.h, C.byref(n)), "sp_batch_last_launches")
        return n.value

    def close(self):
        if self.h:
            lib().sp_batch_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def info_array(info) -> np.ndarray:
    """sp_solve_info[] -> structured numpy view (status, outer, inner, relres)."""
    return np.array([(i.status, i.outer_its, i.inner_its, i.relres) for i in info],
                    dtype=[("status", "i4"), ("outer", "i4"), ("inner", "i4"), ("relres", "f8")])


# ------------------------------------------------------------------ serving

def server_opts(**kw) -> sp_server_opts:
    o = sp_server_opts()
    lib().sp_server_opts_default(C.byref(o))
    names = {f[0] for f in sp_server_opts._fields_}
    for k, v in kw.items():
        if k not in names:
            raise TypeError(f"unknown server option {k!r}")
        setattr(o, k, v)
    return o


class Server:
    """Device-resident request loop over resident RVE geometries."""

    def __init__(self, descs, **opts):
        self.n = len(descs)
        self.descs = (sp_rve_desc * self.n)(*descs)
        self.opts = server_opts(**opts)
        self.h = _vp()
        check(lib().sp_server_create(self.n, self.descs, C.byref(self.opts), C.byref(self.h)),
              "sp_server_create")

    def start(self):
        check(lib().sp_server_start(self.h), "sp_server_start")

    def submit(self, geometry: int, strain) -> int:
        s = np.ascontiguousarray(strain, dtype=np.float64)
        t = C.c_longlong()
        check(lib().sp_server_submit(self.h, geometry, ptr(s), C.byref(t)), "sp_server_submit")
        return t.value

    def poll(self, ticket: int):
        """(stress[6], tangent[6,6], info) or None while pending."""
        st = np.zeros(6)
        tg = np.zeros(36)
        info = sp_solve_info()
        rc = lib().sp_server_poll(self.h, ticket, ptr(st), ptr(tg), C.byref(info))
        if rc == SP_PENDING:
            return None
        check(rc, "sp_server_poll")
        return st, tg.reshape(6, 6), info

    def wait(self, ticket: int, timeout: float = 60.0):
        import time
        t0 = time.time()
        while True:
            r = self.poll(ticket)
            if r is not None:
                return r
            if time.time() - t0 > timeout:
                raise SputnikError(SP_ERR_TIMEOUT, f"ticket {ticket} not done after {timeout}s")
            time.sleep(1e-4)

    def replay(self, geom, strain, t_arrival, timeout=600.0):
        n = len(geom)
        g = np.ascontiguousarray(geom, dtype=np.int32)
        s = np.ascontiguousarray(strain, dtype=np.float64)
        ta = np.ascontiguousarray(t_arrival, dtype=np.float64)
        td = np.zeros(n)
        st = np.zeros((n, 6))
        tg = np.zeros((n, 36))
        info = (sp_solve_info * n)()
        check(lib().sp_server_replay(self.h, n, ptr(g, _ip), ptr(s), ptr(ta), ptr(td), ptr(st),
                                     ptr(tg), info, timeout), "sp_server_replay")
        return td, st, tg.reshape(n, 6, 6), info

    def status(self):
        """(loop on the device now, launches of the loop so far, requests submitted)."""
        on, n, sub = C.c_int(), C.c_longlong(), C.c_longlong()
        check(lib().sp_server_status(self.h, C.byref(on), C.byref(n), C.byref(sub)),
              "sp_server_status")
        return bool(on.value), n.value, sub.value

    def stop(self):
        check(lib().sp_server_stop(self.h), "sp_server_stop")

    def close(self):
        if self.h:
            lib().sp_server_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------- FE2

class Fe2:
    """FE2 cantilever step (sp_fe2_*): macro Newton loop on the GPU, micro
    RVEs through the serving loop."""

    def __init__(self, rves, gp_rve=None, **kw):
        self.d = sp_fe2_desc()
        lib().sp_fe2_desc_default(C.byref(self.d))
        names = {f[0] for f in sp_fe2_desc._fields_}
        for k, v in kw.items():
            if k not in names or k in ("rves", "gp_rve", "nrve"):
                raise TypeError(f"unknown FE2 option {k!r}")
            if k in ("n", "len", "traction"):
                getattr(self.d, k)[:] = v
            else:
                setattr(self.d, k, v)
        self._rves = (sp_rve_desc * len(rves))(*rves)
        self.d.nrve = len(rves)
        self.d.rves = self._rves
        self._gp = None
        if gp_rve is not None:
            self._gp = np.ascontiguousarray(gp_rve, dtype=np.int32)
            self.d.gp_rve = self._gp.ctypes.data_as(C.POINTER(C.c_int))
        self.h = _vp()
        check(lib().sp_fe2_create(C.byref(self.d), C.byref(self.h)), "sp_fe2_create")
        n = list(self.d.n)
        self.ndof = 3 * (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
        self.ngp = 8 * n[0] * n[1] * n[2]

    def run(self) -> sp_fe2_info:
        info = sp_fe2_info()
        check(lib().sp_fe2_run(self.h, C.byref(info)), "sp_fe2_run")
        return info

    def displacement(self) -> np.ndarray:
        u = np.zeros(self.ndof)
        check(lib().sp_fe2_displacement(self.h, ptr(u)), "sp_fe2_displacement")
        return u

    def gp_rve(self) -> np.ndarray:
        g = np.zeros(self.ngp, dtype=np.int32)
        check(lib().sp_fe2_gp_rve(self.h, ptr(g, _ip)), "sp_fe2_gp_rve")
        return g

    def micro_tangents(self) -> np.ndarray:
        Cm = np.zeros((self.d.nrve, 6, 6))
        check(lib().sp_fe2_micro_tangents(self.h, ptr(Cm)), "sp_fe2_micro_tangents")
        return Cm

    def close(self):
        if self.h:
            lib().sp_fe2_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

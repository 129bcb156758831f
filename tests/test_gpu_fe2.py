"""The FE2 step (sp_fe2_*): the GPU macro Newton loop against the CPU FE2
oracle (oracle/fe2.py) fed with the oracle's own micro tangents, and the
per-Gauss-point serving mode against the linear-micro mode."""
import ctypes as C

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import fe2 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, LEN, TRAC = (6, 2, 2), (3.0, 1.0, 1.0), (0.0, 0.0, -1e6)


def rves():
    rng = np.random.default_rng(11)
    out = []
    for n in (3, 4, 3):
        ratio = float(np.exp(rng.uniform(np.log(2), np.log(100))))
        out.append(mb.rve_desc(n, float(rng.uniform(0.15, 0.3)), (1e9, 1e9 * ratio),
                               (float(rng.uniform(0.2, 0.35)), float(rng.uniform(0.2, 0.35)))))
    return out


def oracle_tangent(d):
    m = O.cube_mesh(d.n[0])
    et = O.fiber_types(m, [1, 1], d.radius)
    Cm, _ = O.fd_tangent(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), np.zeros(6), rtol=1e-12,
                         lin_rtol=1e-13)
    return Cm


def gp_binding():
    return np.random.default_rng(5).integers(0, 3, size=8 * np.prod(N)).astype(np.int32)


@pytest.mark.parametrize("clip", [1e-6, 0.0])
def test_fe2_linear_matches_oracle(clip):
    R = rves()
    gp = gp_binding()
    f = mb.Fe2(R, gp_rve=gp, n=N, len=LEN, traction=TRAC, newton_its=3, lin_rtol=1e-12,
               strain_clip=clip)
    info = f.run()
    u = f.displacement()
    Cg = f.micro_tangents()
    assert np.array_equal(f.gp_rve(), gp)
    f.close()
    Co = np.array([oracle_tangent(d) for d in R])
    assert np.abs(Cg - Co).max() <= 1e-7 * np.abs(Co).max()
    # the macro loop on the GPU's micro tangents: displacement to 1e-8
    C_gp = Cg[gp].reshape(np.prod(N), 8, 6, 6)
    uo, norms = F.fe2_cantilever(N, LEN, TRAC, C_gp, newton_its=3, strain_clip=clip)
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    assert info.newton_its == 3
    assert abs(info.bnorm[0] - norms[0]) <= 1e-12 * norms[0]
    assert all(info.pcg_its[i] > 0 for i in range(3))
    assert info.micro_requests == len(R)
    # and on the oracle's own tangents: the tangent difference bounds the gap
    uo2, _ = F.fe2_cantilever(N, LEN, TRAC, Co[gp].reshape(np.prod(N), 8, 6, 6), newton_its=3,
                              strain_clip=clip)
    assert np.linalg.norm(u - uo2) <= 1e-6 * np.linalg.norm(uo2)


def test_fe2_per_gauss_point_serving_matches_linear():
    R = rves()
    gp = gp_binding()
    a = mb.Fe2(R, gp_rve=gp, n=N, len=LEN, traction=TRAC, newton_its=2, lin_rtol=1e-12)
    ia = a.run()
    ua = a.displacement()
    a.close()
    b = mb.Fe2(R, gp_rve=gp, n=N, len=LEN, traction=TRAC, newton_its=2, lin_rtol=1e-12,
               micro=mb.SP_FE2_PER_GP)
    ib = b.run()
    ub = b.displacement()
    b.close()
    assert ib.micro_requests == 2 * 8 * np.prod(N)
    assert np.linalg.norm(ua - ub) <= 1e-7 * np.linalg.norm(ua)
    assert abs(ia.tip[2] - ib.tip[2]) <= 1e-7 * abs(ia.tip[2])


def test_fe2_rejects_bad_binding_and_options():
    R = rves()
    d = mb.sp_fe2_desc()
    mb.lib().sp_fe2_desc_default(C.byref(d))
    d.n[:] = N
    d.len[:] = LEN
    arr = (mb.sp_rve_desc * 3)(*R)
    d.nrve, d.rves = 3, arr
    bad = np.full(8 * np.prod(N), 7, dtype=np.int32)
    d.gp_rve = bad.ctypes.data_as(C.POINTER(C.c_int))
    h = mb._vp()
    assert mb.lib().sp_fe2_create(C.byref(d), C.byref(h)) == mb.SP_ERR_RANGE
    d.gp_rve = None
    d.newton_its = 0
    assert mb.lib().sp_fe2_create(C.byref(d), C.byref(h)) == mb.SP_ERR_ARG

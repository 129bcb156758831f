"""Parity at the benchmark workloads' own mesh sizes, GPU against the FP64
oracle (oracle solves at relative residual 1e-12):

  - batched mixed-precision tangent (4096-RVE mix, n in {8,12,16,20}): RVEs of
    n = 16 and n = 20 drawn as in that mix, stencil and assembled operators,
    mixed and FP64 precision;
  - homogenized tangent of one 24^3 RVE (46,875 dof, 6 unit-strain load
    cases), plain one-RVE path and batch, against the oracle's
    homog_calculate_c_tangent restatement (micro/src/homogenize.c:59-94);
  - serving requests on resident geometries of n = 20 and n = 32 against the
    oracle's finite-difference tangent, stencil and assembled operators;
  - periodic conditions on RVEs of n = 12 and n = 16 against the periodic
    oracle;
  - the FE2 step on the 40x10x10 macro cantilever with 64 RVEs of n = 16:
    micro tangents against the oracle, macro displacement against the FE2
    oracle (oracle/fe2.py) on the same tangents.

Tolerances are the suite's: stress and tangent from unit strains within
1e-8 of max|.|, the FD tangent within 1e-7 (the difference quotient
amplifies the 1e-8 residual), displacements within 1e-8 in the 2-norm."""
import numpy as np
import pytest

import madmax_b200 as mb
from oracle import fe2 as F
from oracle import oracle as O
from oracle import periodic as PER
from oracle import pool as OP

pytestmark = pytest.mark.gpu


def mix_rves(seed, sizes):
    """RVEs drawn as in the batched mix: radius U(0.1, 0.35), fibre/matrix
    stiffness ratio log-uniform in [2, 100], Poisson ratios U(0.2, 0.35)."""
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        ratio = float(np.exp(rng.uniform(np.log(2.0), np.log(100.0))))
        out.append(mb.rve_desc(int(n), float(rng.uniform(0.1, 0.35)), (1e9, 1e9 * ratio),
                               (float(rng.uniform(0.2, 0.35)), float(rng.uniform(0.2, 0.35)))))
    return out


def item(d, *extra):
    return (d.n[0], d.radius, (d.E[0], d.E[1]), (d.nu[0], d.nu[1])) + extra


_cache = {}


def oracle_unit_stress(descs):
    """Oracle stress of the 6 unit strains per RVE (cached per RVE)."""
    todo = [d for d in descs if item(d) not in _cache]
    if todo:
        res = OP.run(OP.homogenize, [item(d, np.eye(6)) for d in todo])
        for d, r in zip(todo, res):
            _cache[item(d)] = r
    return [_cache[item(d)] for d in descs]


HEADLINE = mix_rves(2024, [16, 20, 16, 20])


@pytest.mark.parametrize("precision,op", [(mb.SP_PREC_MIXED, mb.SP_OP_STENCIL),
                                          (mb.SP_PREC_FP64, mb.SP_OP_STENCIL),
                                          (mb.SP_PREC_MIXED, mb.SP_OP_ELL)])
def test_batch_n16_n20_match_oracle(precision, op):
    """The sizes that hold most of the batched mix's time, in the batch's
    default CTA shape, every RVE within 1e-8 of the oracle."""
    st_o = oracle_unit_stress(HEADLINE)
    b = mb.Batch(HEADLINE, precision=precision, op=op)
    stress, strain, info = b.homogenize()
    b.close()
    inf = mb.info_array(info)
    assert (inf["status"] == 0).all() and (inf["relres"] <= 1e-8).all(), inf
    for i in range(len(HEADLINE)):
        err = np.abs(stress[i] - st_o[i]).max() / np.abs(st_o[i]).max()
        assert err <= 1e-8, (i, HEADLINE[i].n[0], err)
        assert np.allclose(strain[i], np.eye(6), atol=1e-12)


def cfg2_rve():
    """One 24^3 RVE, fibre radius U(0.15, 0.35) from a seed, matrix E 1e9
    nu 0.3, fibre E 1e10 nu 0.2."""
    rng = np.random.default_rng(24)
    return mb.rve_desc(24, float(rng.uniform(0.15, 0.35)), (1e9, 1e10), (0.3, 0.2))


def test_n24_tangent_plain_and_batch_match_oracle():
    d = cfg2_rve()
    Co = OP.run(OP.unit_tangent, [item(d)])[0]
    r = mb.Rve(d)
    assert r.ndof == 46875
    Cp, ip = r.tangent(rtol=1e-8)
    r.close()
    assert ip.status == 0 and ip.relres <= 1e-8
    assert np.abs(Cp - Co).max() <= 1e-8 * np.abs(Co).max()
    b = mb.Batch([d])
    s, _, info = b.homogenize()
    b.close()
    assert mb.info_array(info)["status"][0] == 0
    # stress of unit strain e_j is column j of the tangent
    assert np.abs(s[0].T - Co).max() <= 1e-8 * np.abs(Co).max()


@pytest.mark.parametrize("op", [mb.SP_OP_STENCIL, mb.SP_OP_ELL])
def test_serving_n20_n32_match_oracle_fd_tangent(op):
    """Resident geometries of n = 20 and n = 32 (107,811 dof), cold and
    warm-started requests, on the stencil and on the assembled operator:
    stress within 1e-8 and FD tangent within 1e-7."""
    G = mix_rves(32, [20, 32])
    s = mb.Server(G, op=op)
    s.start()
    rng = np.random.default_rng(4)
    reqs = [(0, rng.normal(0, 1e-3, 6)), (1, rng.normal(0, 1e-3, 6)),
            (0, rng.normal(0, 1e-3, 6)), (1, rng.normal(0, 1e-3, 6))]
    tickets = [s.submit(g, e) for g, e in reqs]
    got = [s.wait(t, timeout=300) for t in tickets]
    s.stop()
    s.close()
    key = tuple((g, tuple(e)) for g, e in reqs)
    if key not in _cache:
        _cache[key] = OP.run(OP.fd_tangent, [item(G[g], e) for g, e in reqs])
    want = _cache[key]
    for (st, tg, info), (s0, Cm), (g, _) in zip(got, want, reqs):
        assert info.status == 0 and info.relres <= 1e-8, g
        assert np.abs(st - s0).max() <= 1e-8 * np.abs(s0).max(), g
        assert np.abs(tg - Cm).max() <= 1e-7 * np.abs(Cm).max(), g


def test_periodic_n12_n16_match_oracle():
    """Periodic (master-slave) conditions on RVEs of the mix's sizes 12 and
    16, mixed precision, against the periodic oracle's direct solve."""
    descs = mix_rves(77, [12, 16])
    b = mb.Batch(descs, bc=mb.SP_BC_PERIODIC)
    stress, strain, info = b.homogenize()
    b.close()
    inf = mb.info_array(info)
    assert (inf["status"] == 0).all() and (inf["relres"] <= 1e-8).all(), inf
    for i, d in enumerate(descs):
        m = O.cube_mesh(d.n[0])
        et = O.fiber_types(m, [1, 1], d.radius)
        _, st, _ = PER.homogenize_periodic(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), np.eye(6))
        assert np.abs(stress[i] - st).max() <= 1e-8 * np.abs(st).max(), (i, d.n[0])
        assert np.allclose(strain[i], np.eye(6), atol=1e-12)


def cfg5_rves():
    """64 RVEs of n = 16, fibre radius U(0.15, 0.3) from a seed, matrix E 1e9
    nu 0.3, fibre E 1e10 nu 0.2 (the FE2 step's micro structures)."""
    rng = np.random.default_rng(5150)
    return [mb.rve_desc(16, float(rng.uniform(0.15, 0.3)), (1e9, 1e10), (0.3, 0.2))
            for _ in range(64)]


def test_fe2_full_size_matches_oracle():
    """40x10x10 macro hex8 cantilever (14,883 dof, 32,000 Gauss points), every
    Gauss point bound to one of 64 RVEs of n = 16, two Newton iterations.
    Micro tangents against the oracle; the macro displacement against the
    FE2 oracle on the GPU's tangents (1e-8) and on the oracle's (1e-6).
    Without the reference's strain clip the linear problem is solved by the
    first Newton step: the second residual is at the macro PCG tolerance."""
    R = cfg5_rves()
    f = mb.Fe2(R, newton_its=2, lin_rtol=1e-12, strain_clip=0.0)
    info = f.run()
    u = f.displacement()
    gp = f.gp_rve()
    Cg = f.micro_tangents()
    f.close()
    assert info.newton_its == 2 and info.micro_requests == 64
    assert info.bnorm[1] <= 1e-9 * info.bnorm[0]
    res = OP.run(OP.fd_tangent, [item(d, np.zeros(6)) for d in R])
    Co = np.array([c for _, c in res])
    assert np.abs(Cg - Co).max() <= 1e-7 * np.abs(Co).max()
    n = (40, 10, 10)
    uo, norms = F.fe2_cantilever(n, (4.0, 1.0, 1.0), (0.0, 0.0, -1e6),
                                 Cg[gp].reshape(np.prod(n), 8, 6, 6), newton_its=2,
                                 strain_clip=0.0)
    assert abs(info.bnorm[0] - norms[0]) <= 1e-12 * norms[0]
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    uo2, _ = F.fe2_cantilever(n, (4.0, 1.0, 1.0), (0.0, 0.0, -1e6),
                              Co[gp].reshape(np.prod(n), 8, 6, 6), newton_its=2, strain_clip=0.0)
    assert np.linalg.norm(u - uo2) <= 1e-6 * np.linalg.norm(uo2)

"""Parity of the batched persistent path (sp_batch_*): every RVE of a mixed
batch against the oracle at the hot path's 1e-8 relative tolerance, in mixed
(FP32 CG + FP64 refinement) and FP64 precision; results independent of the
batch an RVE is solved in."""
import ctypes as C

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_descs(seed, sizes):
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        Em = 1e9
        ratio = float(np.exp(rng.uniform(np.log(2), np.log(100))))
        out.append(mb.rve_desc(int(n), float(rng.uniform(0.1, 0.35)), (Em, Em * ratio),
                               (float(rng.uniform(0.2, 0.35)), float(rng.uniform(0.2, 0.35)))))
    return out


def oracle_stress(d, strains):
    n = d.n[0]
    m = O.cube_mesh(n)
    et = O.fiber_types(m, [1, 1], d.radius)
    _, st, _, _ = O.homogenize(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), strains,
                               rtol=1e-12, lin_rtol=1e-13)
    return st


@pytest.mark.parametrize("op", [mb.SP_OP_STENCIL, mb.SP_OP_ELL])
@pytest.mark.parametrize("precision", [mb.SP_PREC_MIXED, mb.SP_PREC_FP64])
def test_batch_unit_tangents_match_oracle(precision, op):
    """Both inner operators: the element-type stencil and the assembled ELL."""
    sizes = [2, 3, 4, 5, 6, 8, 3, 7, 4, 6, 5, 2]
    descs = make_descs(42, sizes)
    b = mb.Batch(descs, precision=precision, op=op)
    stress, strain, info = b.homogenize()
    inf = mb.info_array(info)
    assert (inf["status"] == 0).all(), inf
    assert (inf["relres"] <= 1e-8).all()
    eye = np.eye(6)
    for i, d in enumerate(descs):
        st = oracle_stress(d, eye)
        assert np.abs(stress[i] - st).max() <= 1e-8 * np.abs(st).max(), i
        assert np.allclose(strain[i], eye, atol=1e-12)


@pytest.mark.parametrize("nrhs", [1, 4, 7, 8])
def test_batch_custom_strains_and_materials(nrhs):
    descs = make_descs(7, [3, 5, 4, 6])
    rng = np.random.default_rng(nrhs)
    strains = rng.normal(0, 1e-3, size=(len(descs), nrhs, 6))
    mats = np.array([[2e9, 0.28, 3e10, 0.22], [1e9, 0.3, 1e9 * 50, 0.3],
                     [5e9, 0.2, 1e10, 0.35], [1e9, 0.33, 1e11, 0.21]])
    b = mb.Batch(descs, nrhs=nrhs)
    stress, _, info = b.homogenize(np.ascontiguousarray(strains), mats)
    assert (mb.info_array(info)["status"] == 0).all()
    for i, d in enumerate(descs):
        d.E[0], d.nu[0], d.E[1], d.nu[1] = mats[i]
        st = oracle_stress(d, strains[i])
        assert np.abs(stress[i] - st).max() <= 1e-8 * np.abs(st).max()


def test_same_result_alone_and_in_mix():
    """At a fixed CTA shape an RVE's result is bit-identical alone and in a
    mix, and from launch to launch."""
    descs = make_descs(3, [6, 2, 8, 4, 6, 3, 5, 7, 2, 4] * 3)
    big = mb.Batch(descs, threads=512, ctas_per_sm=1)
    s_mix, _, _ = big.homogenize()
    for i in (0, 7, 19):
        alone = mb.Batch([descs[i]], threads=512, ctas_per_sm=1)
        s1, _, _ = alone.homogenize()
        assert np.array_equal(s1[0], s_mix[i])
    # and repeatable launch to launch
    s_again, _, _ = big.homogenize()
    assert np.array_equal(s_again, s_mix)


@pytest.mark.parametrize("threads,ctas,cluster,op", [
    (512, 1, 1, mb.SP_OP_ELL), (512, 2, 1, mb.SP_OP_ELL), (256, 2, 1, mb.SP_OP_ELL),
    (256, 4, 1, mb.SP_OP_ELL), (512, 2, 2, mb.SP_OP_ELL), (512, 1, 4, mb.SP_OP_ELL),
    (512, 2, 8, mb.SP_OP_ELL), (512, 1, 1, mb.SP_OP_STENCIL), (512, 2, 1, mb.SP_OP_STENCIL),
    (256, 2, 1, mb.SP_OP_STENCIL), (256, 4, 1, mb.SP_OP_STENCIL), (1024, 1, 1, mb.SP_OP_STENCIL)])
def test_cta_shapes_agree(threads, ctas, cluster, op):
    """Every CTA shape, and RVEs split over thread-block clusters of 2, 4
    and 8 CTAs, give the oracle's result."""
    descs = make_descs(9, [5, 3, 6, 2, 8, 12])
    b = mb.Batch(descs, threads=threads, ctas_per_sm=ctas, cluster=cluster, op=op)
    s, _, info = b.homogenize()
    assert (mb.info_array(info)["status"] == 0).all()
    for i, d in enumerate(descs):
        st = oracle_stress(d, np.eye(6))
        assert np.abs(s[i] - st).max() <= 1e-8 * np.abs(st).max()


def test_cluster_result_is_deterministic():
    descs = make_descs(21, [6, 10, 4])
    a, _, _ = mb.Batch(descs, cluster=4, op=mb.SP_OP_ELL).homogenize()
    b, _, _ = mb.Batch(descs, cluster=4, op=mb.SP_OP_ELL).homogenize()
    c, _, _ = mb.Batch(descs[1:2], cluster=4, op=mb.SP_OP_ELL).homogenize()
    assert np.array_equal(a, b)
    assert np.array_equal(a[1], c[0])


def test_stencil_and_assembled_agree_on_boxes():
    """Non-cubic meshes (nx != ny != nz, unequal edge lengths): the stencil
    operator and the assembled ELL operator reach the same tangent."""
    descs = make_descs(5, [4, 6, 5, 3])
    for d, n, ln in zip(descs, [(3, 5, 4), (6, 2, 7), (5, 5, 9), (2, 3, 2)],
                        [(1.0, 1.5, 0.8), (2.0, 1.0, 1.0), (1.0, 1.0, 1.7), (0.5, 1.0, 1.0)]):
        d.n[0], d.n[1], d.n[2] = n
        d.len[0], d.len[1], d.len[2] = ln
    a, _, ia = mb.Batch(descs, op=mb.SP_OP_STENCIL).homogenize()
    b, _, ib = mb.Batch(descs, op=mb.SP_OP_ELL).homogenize()
    assert (mb.info_array(ia)["status"] == 0).all() and (mb.info_array(ib)["status"] == 0).all()
    for i in range(len(descs)):
        assert np.abs(a[i] - b[i]).max() <= 2e-8 * np.abs(b[i]).max(), i


def test_unknown_batch_option_is_rejected():
    with pytest.raises(TypeError):
        mb.batch_opts(oprator=1)


# ------------------------------------------------- periodic conditions ---

from oracle import periodic as PER  # noqa: E402


def test_periodic_tangents_match_oracle():
    """Periodic (master-slave) conditions on the stencil path against the
    CPU periodic oracle at 1e-8, in both precisions."""
    descs = make_descs(31, [2, 3, 4, 5, 6, 8, 4])
    for prec in (mb.SP_PREC_MIXED, mb.SP_PREC_FP64):
        s, strain, info = mb.Batch(descs, bc=mb.SP_BC_PERIODIC, precision=prec).homogenize()
        inf = mb.info_array(info)
        assert (inf["status"] == 0).all() and (inf["relres"] <= 1e-8).all()
        for i, d in enumerate(descs):
            m = O.cube_mesh(d.n[0])
            et = O.fiber_types(m, [1, 1], d.radius)
            _, st, _ = PER.homogenize_periodic(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]),
                                               np.eye(6))
            assert np.abs(s[i] - st).max() <= 1e-8 * np.abs(st).max(), (prec, i)
            assert np.allclose(strain[i], np.eye(6), atol=1e-12)


def test_periodic_homogeneous_box_gives_D():
    """A homogeneous RVE (both materials equal) under periodic conditions is
    a patch test: the fluctuation vanishes and <sigma> = D eps exactly, on
    non-cubic boxes too."""
    descs = make_descs(3, [3, 4, 5])
    for d, n, ln in zip(descs, [(3, 4, 2), (4, 4, 4), (6, 2, 3)],
                        [(1.0, 1.3, 0.7), (1.0, 1.0, 1.0), (2.0, 0.5, 1.0)]):
        d.n[0], d.n[1], d.n[2] = n
        d.len[0], d.len[1], d.len[2] = ln
        d.E[1], d.nu[1] = d.E[0], d.nu[0]
    s, _, info = mb.Batch(descs, bc=mb.SP_BC_PERIODIC).homogenize()
    assert (mb.info_array(info)["status"] == 0).all()
    for i, d in enumerate(descs):
        D = np.zeros(36)
        O.lib().orc_iso_D(3, d.E[0], d.nu[0], O.ptr(D))
        assert np.abs(s[i] - D.reshape(6, 6)).max() <= 1e-9 * d.E[0], i


def test_periodic_is_softer_than_affine():
    """Hill bounds: C_affine - C_periodic is positive semi-definite."""
    descs = make_descs(8, [6, 8])
    sa, _, _ = mb.Batch(descs).homogenize()
    sp, _, _ = mb.Batch(descs, bc=mb.SP_BC_PERIODIC).homogenize()
    for i in range(len(descs)):
        dC = sa[i].T - sp[i].T
        ev = np.linalg.eigvalsh((dC + dC.T) / 2)
        assert ev.min() >= -1e-7 * np.abs(sa[i]).max()
        assert ev.max() > 1e-3 * np.abs(sa[i]).max()


def test_periodic_rejects_assembled_operator_and_thin_meshes():
    import ctypes as C
    descs = make_descs(1, [4])
    arr = (mb.sp_rve_desc * 1)(*descs)
    h = mb._vp()
    o = mb.batch_opts(bc=mb.SP_BC_PERIODIC, op=mb.SP_OP_ELL)
    assert mb.lib().sp_batch_create(1, arr, C.byref(o), C.byref(h)) == mb.SP_ERR_ARG
    descs[0].n[2] = 1
    arr = (mb.sp_rve_desc * 1)(*descs)
    o = mb.batch_opts(bc=mb.SP_BC_PERIODIC)
    assert mb.lib().sp_batch_create(1, arr, C.byref(o), C.byref(h)) == mb.SP_ERR_ARG


def test_default_shape_per_operator():
    """The fixed defaults, when the autotuner is off: 512 x 1 for the stencil
    (128 registers a thread), 512 x 2 for the assembled operator."""
    descs = make_descs(2, [4, 5])
    off = mb.SP_TUNE_OFF
    assert mb.Batch(descs, tune=off).shape()[:2] == (512, 1)
    assert mb.Batch(descs, op=mb.SP_OP_ELL, tune=off).shape()[:2] == (512, 2)
    assert mb.Batch(descs, bc=mb.SP_BC_PERIODIC, tune=off).shape()[:2] == (512, 1)
    assert mb.Batch(descs, precision=mb.SP_PREC_FP64, tune=off).shape()[:2] == (512, 1)
    assert mb.Batch(descs, op=mb.SP_OP_ELL, precision=mb.SP_PREC_FP64,
                    tune=off).shape()[:2] == (512, 2)
    assert mb.lib().sp_batch_create(2, (mb.sp_rve_desc * 2)(*descs),
                                    C.byref(mb.batch_opts(tune=5)),
                                    C.byref(mb._vp())) == mb.SP_ERR_ARG


# --------------------------------------------------- edge and full sizes ---

def test_single_element_and_thin_meshes():
    """n = 1 (every node on the boundary: nothing to solve) and meshes one
    element thick agree with the oracle; an empty batch is refused."""
    import ctypes as C
    descs = make_descs(12, [1, 2, 1])
    descs[1].n[0], descs[1].n[1], descs[1].n[2] = 1, 3, 2
    s, strain, info = mb.Batch(descs).homogenize()
    inf = mb.info_array(info)
    assert (inf["status"] == 0).all() and (inf["inner"][[0, 2]] == 0).all()
    for i in (0, 2):
        d = descs[i]
        m = O.cube_mesh(1)
        et = O.fiber_types(m, [1, 1], d.radius)
        _, st, _, _ = O.homogenize(m, et, (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), np.eye(6),
                                   rtol=1e-12, lin_rtol=1e-13)
        assert np.abs(s[i] - st).max() <= 1e-8 * np.abs(st).max()
    e, _, _ = mb.Batch([descs[1]], op=mb.SP_OP_ELL).homogenize()
    assert np.abs(s[1] - e[0]).max() <= 2e-8 * np.abs(e[0]).max()
    h = mb._vp()
    arr = (mb.sp_rve_desc * 1)(*descs[:1])
    assert mb.lib().sp_batch_create(0, arr, None, C.byref(h)) == mb.SP_ERR_ARG


def test_large_rve_size_independent_properties():
    """A 40^3 RVE (206,763 dof), too large for the CPU oracle in a test:
    the stencil and assembled operators agree, the tangent is symmetric
    (major symmetry of the homogenized stiffness), its diagonal is positive,
    and the periodic tangent is bounded by it (Hill).  The two operators are
    compared at a 1e-10 residual: at 1e-8 the tangents of two different FP32
    iterations of this large RVE can differ by ~1e-7 of their scale."""
    d = make_descs(40, [40])[0]
    a, _, ia = mb.Batch([d], rtol=1e-10).homogenize()
    b, _, ib = mb.Batch([d], op=mb.SP_OP_ELL, rtol=1e-10).homogenize()
    p, _, ip = mb.Batch([d], bc=mb.SP_BC_PERIODIC).homogenize()
    for inf in (ia, ib, ip):
        assert (mb.info_array(inf)["status"] == 0).all()
    Ca, Cb, Cp = a[0].T, b[0].T, p[0].T
    scale = np.abs(Ca).max()
    assert np.abs(Ca - Cb).max() <= 2e-8 * scale
    assert np.abs(Ca - Ca.T).max() <= 1e-7 * scale
    assert (np.diag(Ca) > 0).all()
    dC = Ca - Cp
    assert np.linalg.eigvalsh((dC + dC.T) / 2).min() >= -1e-7 * scale


def test_larger_sizes_stencil_agrees_with_assembled():
    """The bench's larger sizes and beyond (n = 16 ... 28) on the stencil at
    both one-CTA-per-SM shapes give the assembled operator's tangent, which
    is tested against the oracle.  Compared at a 1e-10 residual, so that the
    two operators' different FP32 iterations cannot separate the tangents by
    more than the tolerance."""
    descs = make_descs(77, [16, 20, 24, 28, 20])
    for threads in (1024, 512):
        a, _, ia = mb.Batch(descs, threads=threads, ctas_per_sm=1, rtol=1e-10).homogenize()
        assert (mb.info_array(ia)["status"] == 0).all()
        if threads == 1024:
            b, _, ib = mb.Batch(descs, op=mb.SP_OP_ELL, rtol=1e-10).homogenize()
            assert (mb.info_array(ib)["status"] == 0).all()
        for i in range(len(descs)):
            assert np.abs(a[i] - b[i]).max() <= 2e-8 * np.abs(b[i]).max(), (threads, i)


def test_voxel_materials_match_oracle():
    """Arbitrary two-material voxel micro-structures (random element
    materials, not invariant along z: every material pattern a node can
    see), set with sp_batch_set_etype: the stencil's pattern tables, the
    assembled operator and FP64 all give the oracle's tangent."""
    rng = np.random.default_rng(17)
    descs = make_descs(23, [3, 4, 5, 6])
    ets = [(rng.random(d.n[0] ** 3) < 0.4).astype(np.uint8) for d in descs]
    for kw in ({}, {"op": mb.SP_OP_ELL}, {"precision": mb.SP_PREC_FP64},
               {"threads": 1024, "ctas_per_sm": 1}):
        b = mb.Batch(descs, **kw)
        for i, et in enumerate(ets):
            b.set_etype(i, et)
        s, _, info = b.homogenize()
        assert (mb.info_array(info)["status"] == 0).all(), kw
        for i, d in enumerate(descs):
            m = O.cube_mesh(d.n[0])
            _, st, _, _ = O.homogenize(m, ets[i], (d.E[0], d.E[1]), (d.nu[0], d.nu[1]), np.eye(6),
                                       rtol=1e-12, lin_rtol=1e-13)
            assert np.abs(s[i] - st).max() <= 1e-8 * np.abs(st).max(), (kw, i)


def test_set_etype_rejects_bad_input():
    b = mb.Batch(make_descs(2, [3]))
    with pytest.raises(mb.SputnikError):
        b.set_etype(1, np.zeros(27, np.uint8))
    with pytest.raises(mb.SputnikError):
        b.set_etype(0, np.full(27, 2, np.uint8))


@pytest.mark.parametrize("op", [mb.SP_OP_STENCIL, mb.SP_OP_ELL])
def test_autotuned_shape_is_measured_cached_and_correct(op):
    """A batch whose shape is left open is timed on every instantiated CTA
    shape; the fastest is launched, the choice is cached for the next batch
    of the same kind, and results match the oracle; a batch whose shape is
    given is not tuned."""
    descs = make_descs(77, [9, 7, 9, 8, 6, 9, 5, 9] * 40)
    a = mb.Batch(descs, op=op)
    rep = a.tune_report()
    assert rep and len(rep["candidates"]) >= 2
    rates = [c["rate"] for c in rep["candidates"]]
    best = rep["candidates"][int(np.argmax(rates))]
    assert rep["chosen"] == {"threads": best["threads"], "ctas_per_sm": best["ctas_per_sm"]}
    t, c, g = a.shape()
    assert (t, c) == (best["threads"], best["ctas_per_sm"]) and g % c == 0
    s, _, info = a.homogenize()
    a.close()
    assert (mb.info_array(info)["status"] == 0).all()
    for i in (0, 1, 4):
        st = oracle_stress(descs[i], np.eye(6))
        assert np.abs(s[i] - st).max() <= 1e-8 * np.abs(st).max()
    b = mb.Batch(descs, op=op)
    rb = b.tune_report()
    b.close()
    assert rb["from_cache"] and rb["chosen"] == rep["chosen"]
    fixed = mb.Batch(descs[:4], op=op, threads=512, ctas_per_sm=2)
    assert fixed.tune_report() == {} and fixed.shape()[:2] == (512, 2)
    fixed.close()
    off = mb.Batch(descs[:4], op=op, tune=mb.SP_TUNE_OFF)
    assert off.tune_report() == {}
    off.close()


def test_batch_launch_captured_in_a_cuda_graph():
    """A batch launch (a counter reset and one persistent kernel on the
    caller's stream) is captured in a CUDA graph and replayed: the replays
    give the same results as a direct launch, bit for bit, and match the
    oracle."""
    import torch
    descs = make_descs(13, [6, 8, 5, 7, 4, 8])
    b = mb.Batch(descs, threads=512, ctas_per_sm=1)
    s = torch.cuda.Stream()
    sp = C.c_void_p(s.cuda_stream)
    direct = np.zeros((len(descs), 6, 6))
    b.launch(sp)
    b.download(direct, None, None, sp)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(sp)
    for _ in range(2):
        out = np.zeros((len(descs), 6, 6))
        info = (mb.sp_solve_info * len(descs))()
        g.replay()
        torch.cuda.synchronize()
        b.download(out, None, info, sp)
        s.synchronize()
        assert (mb.info_array(info)["status"] == 0).all()
        assert np.array_equal(out, direct)
    del g
    b.close()
    for i in (0, 3):
        st = oracle_stress(descs[i], np.eye(6))
        assert np.abs(direct[i] - st).max() <= 1e-8 * np.abs(st).max()
